"""Seeded synthetic case generators (geometry, boundary records, initial state).

There is no public dataset for this path: the reference's own test cases define the shapes
(test/1D/Sod79, test/1D/ShuOsher-LIMO3, test/2D/euler/{ramp-channel, chang-nozzle,
planar-nozzle}); these generators build cases with those layouts and the workload sizes of
the benchmark configurations, seeded with numpy's PCG64 at stated seeds.

Array conventions (C order, matching the Fortran memory order of the reference arrays):
  nodes: (nj+1, ni+1, 2)  == node(2, 0:ni, 0:nj)
  area:  (nj+1, ni+1)     == Cross_Section(0:ni, 0:nj)
  prim:  (nj, ni, 4)      interior cells, variables rho, u, v, p
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ._abi import NORMAL_DIR

BASE_SEED = 20261203


@dataclass
class BlockSpec:
    ni: int
    nj: int
    nodes: np.ndarray
    prim: np.ndarray
    area: Optional[np.ndarray] = None

    def prim_ghost(self, ghosts: Optional[float] = 0.0) -> np.ndarray:
        """The interior state embedded in the reference layout P(4, -1:ni+2, -1:nj+2); the ghost
        layers hold `ghosts` (None leaves them unset: the C ABI never reads them)."""
        P = np.empty((self.nj + 4, self.ni + 4, 4)) if ghosts is None else \
            np.full((self.nj + 4, self.ni + 4, 4), ghosts)
        P[2:self.nj + 2, 2:self.ni + 2, :] = self.prim
        return P

    @property
    def cells(self) -> int:
        return self.ni * self.nj


@dataclass
class CaseSpec:
    name: str
    blocks: list
    bcs: list
    options: dict = field(default_factory=dict)
    meta: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return sum(b.cells for b in self.blocks)


# ------------------------------------------------------------------------------------------
# boundary-record helpers (bc.txt layout: header b,i,j,f,type + property fields)
# ------------------------------------------------------------------------------------------
def edge_records(b: int, ni: int, nj: int, faces: dict) -> list:
    """Records for the 4 edges of block b in bc.txt order (face 1..4). faces[f] is
    (type, props) or a callable (k) -> (type, props) for per-cell types."""
    recs = []
    for f in (1, 2, 3, 4):
        if f not in faces:
            continue
        n = nj if f <= 2 else ni
        for k in range(1, n + 1):
            spec = faces[f](k) if callable(faces[f]) else faces[f]
            typ, props = spec
            if f == 1:
                i, j = 1, k
            elif f == 2:
                i, j = ni, k
            elif f == 3:
                i, j = k, 1
            else:
                i, j = k, nj
            r = {"b": b, "i": i, "j": j, "f": f, "type": typ}
            r.update(props)
            recs.append(r)
    return recs


def stagnation_props(T0: float, p0: float) -> dict:
    return {"T0": T0, "p0": p0, "alpha": NORMAL_DIR, "rel_fac": 1.0}


def supersonic_props(mach: float, T: float, p: float) -> dict:
    return {"mach": mach, "T0": T, "pamb": p, "alpha": NORMAL_DIR, "rel_fac": 1.0}


# ------------------------------------------------------------------------------------------
# quasi-1D isentropic flow, used for nozzle initial states
# ------------------------------------------------------------------------------------------
def area_mach(M, g):
    return (1.0 / M) * ((2.0 / (g + 1)) * (1.0 + 0.5 * (g - 1) * M * M)) ** ((g + 1) / (2 * (g - 1)))


def mach_of_area(ar: np.ndarray, supersonic: np.ndarray, g: float) -> np.ndarray:
    ar = np.maximum(np.asarray(ar, dtype=float), 1.0)
    lo = np.where(supersonic, 1.0 + 1e-9, 1e-7)
    hi = np.where(supersonic, 80.0, 1.0 - 1e-9)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        f = area_mach(mid, g) - ar
        # area ratio decreases with M below 1 and increases above 1
        go_up = np.where(supersonic, f < 0, f > 0)
        lo = np.where(go_up, mid, lo)
        hi = np.where(go_up, hi, mid)
    return 0.5 * (lo + hi)


def isentropic_state(M, p0, T0, R, g):
    tf = 1.0 + 0.5 * (g - 1) * M * M
    T = T0 / tf
    p = p0 * tf ** (-g / (g - 1))
    rho = p / (R * T)
    u = M * np.sqrt(g * R * T)
    return rho, u, p


# ------------------------------------------------------------------------------------------
# configurations
# ------------------------------------------------------------------------------------------
def riemann_1d(ni: int = 1024, nj: int = 4, seed: int = BASE_SEED, states=None,
               limiter: str = "minmod", t_end: float = 0.15) -> CaseSpec:
    """1-D Riemann problem on a ni x nj planar block, x in [0,1], y in [0, nj/ni] (square
    cells), diaphragm at x = 0.5; BC 400 on the i ends, 300 on the j sides
    (test/1D/Sod79 layout). rho_L, p_L ~ U[0.5, 2]; rho_R, p_R ~ U[0.05, 0.5]; u = v = 0."""
    rng = np.random.default_rng(seed)
    if states is None:
        rl, pl = rng.uniform(0.5, 2.0, 2)
        rr, pr = rng.uniform(0.05, 0.5, 2)
    else:
        rl, pl, rr, pr = states
    xn = np.linspace(0.0, 1.0, ni + 1)
    yn = np.linspace(0.0, nj / ni, nj + 1)
    nodes = np.stack(np.meshgrid(xn, yn), axis=-1)
    xc = 0.5 * (xn[:-1] + xn[1:])
    prim = np.zeros((nj, ni, 4))
    left = xc < 0.5
    prim[:, :, 0] = np.where(left, rl, rr)
    prim[:, :, 3] = np.where(left, pl, pr)
    blk = BlockSpec(ni, nj, nodes, prim)
    bcs = edge_records(1, ni, nj, {1: (400, {}), 2: (400, {}), 3: (300, {}), 4: (300, {})})
    opts = dict(limiter=limiter, riemann="HLLC", n_rk=3, cfl=0.5, time_accurate=1,
                time_threshold=t_end, gas_R=287.0, gas_gamma=1.4)
    return CaseSpec("riemann1d", [blk], bcs, opts,
                    {"states": (rl, 0.0, pl, rr, 0.0, pr), "x0": 0.5, "t_end": t_end})


def shuosher(ni: int = 400, runiv: float = 8314.46, gamma: float = 1.4) -> CaseSpec:
    """Shu-Osher problem with the layout of test/1D/ShuOsher-LIMO3/gen_case.py:19-35,47-53
    (x in [-5,5], 1 cell row, BC 400 on the i ends and 300 on the j sides) and the constant-cp
    Air table of test/common/Air (cp = 1004.5, W = 28.970418). The reference binary's outputs
    are reproduced with gamma = 1.4 exactly (the table's cp/(cp-R) = 1.399996 fits them 1000x
    worse), so gamma defaults to 1.4; R only scales T, which cancels in the closure."""
    nj = 1
    xn = np.array([-5.0 + i * (10.0 / ni) for i in range(ni + 1)])
    yn = np.array([0.0, 1.0])
    nodes = np.stack(np.meshgrid(xn, yn), axis=-1)
    xc = 0.5 * (xn[:-1] + xn[1:])
    prim = np.zeros((nj, ni, 4))
    post = xc < -4.0
    prim[0, :, 0] = np.where(post, 3.857143, 1.0 + 0.2 * np.sin(5.0 * xc))
    prim[0, :, 1] = np.where(post, 2.629369, 0.0)
    prim[0, :, 3] = np.where(post, 10.33333, 1.0)
    R = runiv / 28.970418
    blk = BlockSpec(ni, nj, nodes, prim)
    bcs = edge_records(1, ni, nj, {1: (400, {}), 2: (400, {}), 3: (300, {}), 4: (300, {})})
    opts = dict(riemann="HLLC", n_rk=3, cfl=0.5, time_accurate=1, time_threshold=1.8,
                gas_R=R, gas_gamma=gamma)
    return CaseSpec("shuosher", [blk], bcs, opts, {"xc": xc})


def ramp(ni: int = 1536, nj: int = 512, seed: int = BASE_SEED + 1, theta_deg=None,
         mach=None, top_bc: int = 400) -> CaseSpec:
    """Supersonic flow over a compression ramp (test/2D/euler/ramp-channel layout: BC 405
    inflow, 400 outflow, 300 lower wall; the upper boundary is 400 unless top_bc says 300).
    Domain length L = 1, height H = 0.5, corner at x = 0.3 L, angle ~ U[5, 15] deg, inflow
    Mach ~ U[2, 3] at T = 300 K, p = 1e5 Pa; gamma = 1.4, R = 287."""
    rng = np.random.default_rng(seed)
    th = math.radians(theta_deg if theta_deg is not None else rng.uniform(5.0, 15.0))
    M = mach if mach is not None else rng.uniform(2.0, 3.0)
    L, H, xc0 = 1.0, 0.5, 0.3
    R, g, T, p = 287.0, 1.4, 300.0, 1.0e5
    xn = np.linspace(0.0, L, ni + 1)
    yw = np.maximum(xn - xc0 * L, 0.0) * math.tan(th)
    eta = np.linspace(0.0, 1.0, nj + 1)
    X = np.broadcast_to(xn[None, :], (nj + 1, ni + 1))
    Y = yw[None, :] + (H - yw[None, :]) * eta[:, None]
    nodes = np.stack([X, Y], axis=-1).copy()
    rho = p / (R * T)
    a = math.sqrt(g * R * T)
    prim = np.zeros((nj, ni, 4))
    prim[..., 0] = rho
    prim[..., 1] = M * a
    prim[..., 3] = p
    blk = BlockSpec(ni, nj, nodes, prim)
    bcs = edge_records(1, ni, nj, {1: (405, supersonic_props(M, T, p)), 2: (400, {}),
                                   3: (300, {}), 4: (top_bc, {})})
    opts = dict(limiter="vanleer", riemann="HLLC", n_rk=3, cfl=0.5, time_accurate=0,
                gas_R=R, gas_gamma=g)
    return CaseSpec("ramp", [blk], bcs, opts, {"theta": th, "mach": M})


def nozzle_axi(ni: int = 512, nj: int = 128, nblocks: int = 4, seed: int = BASE_SEED + 2,
               p0=None, T0=None) -> CaseSpec:
    """Axisymmetric converging-diverging nozzle, wall radius r(x) = 1 + 1.5 (x-1)^2 on
    x in [0,3], throat at x = 1, split in x into nblocks blocks stitched by BC 101
    (test/2D/euler/chang-nozzle layout: 401 inflow, 400 outflow, 300 axis and wall).
    p0 ~ U[2, 10] bar, T0 ~ U[300, 800] K; quasi-1D isentropic initial state with the flow
    angle interpolated linearly from the axis (0) to the wall slope."""
    rng = np.random.default_rng(seed)
    p0 = p0 if p0 is not None else rng.uniform(2e5, 10e5)
    T0 = T0 if T0 is not None else rng.uniform(300.0, 800.0)
    R, g = 287.0, 1.4
    blocks, bcs = [], []
    xs = np.linspace(0.0, 3.0, nblocks + 1)
    for k in range(nblocks):
        xn = np.linspace(xs[k], xs[k + 1], ni + 1)
        rw = 1.0 + 1.5 * (xn - 1.0) ** 2
        eta = np.linspace(0.0, 1.0, nj + 1)
        X = np.broadcast_to(xn[None, :], (nj + 1, ni + 1))
        Y = rw[None, :] * eta[:, None]
        nodes = np.stack([X, Y], axis=-1).copy()
        xc = 0.5 * (xn[:-1] + xn[1:])
        ar = (1.0 + 1.5 * (xc - 1.0) ** 2) ** 2
        M = mach_of_area(ar, xc > 1.0, g)
        rho, q, p = isentropic_state(M, p0, T0, R, g)
        # flow direction interpolated between the axis (0) and the wall slope dr/dx
        yc = 0.25 * (Y[:-1, :-1] + Y[1:, :-1] + Y[:-1, 1:] + Y[1:, 1:])
        rc = 1.0 + 1.5 * (xc - 1.0) ** 2
        ang = np.arctan(3.0 * (xc - 1.0))[None, :] * (yc / rc[None, :])
        prim = np.zeros((nj, ni, 4))
        prim[..., 0] = rho[None, :]
        prim[..., 1] = q[None, :] * np.cos(ang)
        prim[..., 2] = q[None, :] * np.sin(ang)
        prim[..., 3] = p[None, :]
        blocks.append(BlockSpec(ni, nj, nodes, prim))
        b = k + 1
        f1 = (401, stagnation_props(T0, p0)) if k == 0 else \
            (lambda kk, b=b: (101, dict(bs=b - 1, is_=ni, js=kk, fs=2, d11=1, d12=0, d21=0, d22=1)))
        f2 = (400, {}) if k == nblocks - 1 else \
            (lambda kk, b=b: (101, dict(bs=b + 1, is_=1, js=kk, fs=1, d11=1, d12=0, d21=0, d22=1)))
        bcs += edge_records(b, ni, nj, {1: f1, 2: f2, 3: (300, {}), 4: (300, {})})
    # The wall opens to 80 degrees at the exit; minmod, CFL 0.3 and a 200-step CFL ramp
    # (cfl-rise-threshold) keep the start-up transient positive.
    opts = dict(limiter="minmod", riemann="HLLC", n_rk=3, cfl=0.3, time_accurate=0, rampa_iter=200,
                source="axisymmetric", res_threshold=1e-10, gas_R=R, gas_gamma=g)
    return CaseSpec("nozzle_axi", blocks, bcs, opts, {"p0": p0, "T0": T0})


def area_nozzle(ni: int, nj: int, k: float, xt: float, p0: float, T0: float) -> CaseSpec:
    """Quasi-2D area-variation nozzle (test/2D/euler/planar-nozzle layout: 401 inflow, 400
    outflow, 300/300 sides, nodal Cross_Section): x in [0,1], y in [0, 0.1],
    A(x) = A_t (1 + k (x - x_t)^2), quasi-1D isentropic initial state."""
    R, g = 287.0, 1.4
    xn = np.linspace(0.0, 1.0, ni + 1)
    yn = np.linspace(0.0, 0.1, nj + 1)
    nodes = np.stack(np.meshgrid(xn, yn), axis=-1)
    area_n = 1.0 + k * (xn - xt) ** 2
    area = np.broadcast_to(area_n[None, :], (nj + 1, ni + 1)).copy()
    xc = 0.5 * (xn[:-1] + xn[1:])
    M = mach_of_area(1.0 + k * (xc - xt) ** 2, xc > xt, g)
    rho, u, p = isentropic_state(M, p0, T0, R, g)
    prim = np.zeros((nj, ni, 4))
    prim[..., 0] = rho[None, :]
    prim[..., 1] = u[None, :]
    prim[..., 3] = p[None, :]
    blk = BlockSpec(ni, nj, nodes, prim, area)
    bcs = edge_records(1, ni, nj, {1: (401, stagnation_props(T0, p0)), 2: (400, {}),
                                   3: (300, {}), 4: (300, {})})
    opts = dict(limiter="vanleer", riemann="HLLC", n_rk=3, cfl=0.5, time_accurate=0,
                source="area_variation", gas_R=R, gas_gamma=g)
    return CaseSpec("area_nozzle", [blk], bcs, opts,
                    {"k": k, "xt": xt, "p0": p0, "T0": T0})


def planar_nozzle_area(x):
    """Cross-section of the reference's planar-nozzle case (test/2D/euler/planar-nozzle/
    gen_case.py:30-35): throat A_t = 1 at x_t = 0.4 on x in [0, 1], inlet A = 2, exit A = 2.5,
    half-cosine blends on each side, so that dA/dx = 0 at the throat."""
    x = np.asarray(x, dtype=np.float64)
    up = 1.0 + (2.0 - 1.0) * 0.5 * (1.0 + np.cos(np.pi * x / 0.4))
    down = 1.0 + (2.5 - 1.0) * 0.5 * (1.0 - np.cos(np.pi * (x - 0.4) / 0.6))
    return np.where(x <= 0.4, up, down)


def planar_nozzle(ni: int = 200, nj: int = 4) -> CaseSpec:
    """The reference's planar-nozzle steady case (test/2D/euler/planar-nozzle/gen_case.py:19-94,
    input.ini): x in [0, 1], y in [0, 0.1], the cross-section above as nodal Cross_Section,
    constant-cp air (c_p = 1004.5, W = 28.970418, Runiv = 8314.462618), stagnation inflow
    p0 = 1e6 Pa, T0 = 300 K (BC 401, 'normal'), extrapolation outflow (400), symmetry sides (300),
    the quasi-1D isentropic state as initial condition (subsonic before the throat, supersonic
    after); van Leer MUSCL + HLLC, SSP-RK3, CFL 0.5 with a 50-iteration ramp, IRS beta 0.5, local
    time steps, area-variation sources, 40000 iterations at most."""
    R = 8314.462618 / 28.970418
    g = 1004.5 / (1004.5 - R)
    p0, T0 = 1.0e6, 300.0
    xn = np.linspace(0.0, 1.0, ni + 1)
    yn = np.linspace(0.0, 0.1, nj + 1)
    nodes = np.stack(np.meshgrid(xn, yn), axis=-1)
    area = np.broadcast_to(planar_nozzle_area(xn)[None, :], (nj + 1, ni + 1)).copy()
    xc = 0.5 * (xn[:-1] + xn[1:])
    M = mach_of_area(planar_nozzle_area(xc), xc > 0.4, g)
    rho, u, p = isentropic_state(M, p0, T0, R, g)
    prim = np.zeros((nj, ni, 4))
    prim[..., 0] = rho[None, :]
    prim[..., 1] = u[None, :]
    prim[..., 3] = p[None, :]
    blk = BlockSpec(ni, nj, nodes, prim, area)
    bcs = edge_records(1, ni, nj, {1: (401, stagnation_props(T0, p0)), 2: (400, {}),
                                   3: (300, {}), 4: (300, {})})
    opts = dict(limiter="vanleer", riemann="HLLC", n_rk=3, cfl=0.5, rampa_iter=50, time_accurate=0,
                irs_beta=0.5, source="area_variation", itermax=40000, gas_R=R, gas_gamma=g)
    return CaseSpec("planar_nozzle", [blk], bcs, opts, {"xc": xc, "p0": p0, "T0": T0})


def area_nozzle_batch(n: int = 4096, seed: int = BASE_SEED + 3, nx_range=(64, 1024),
                      ny_range=(8, 64)) -> list:
    """The batched workload: n independent area-variation nozzles with
    Nx = clip(round(exp(N(ln 256, 0.6))), 64, 1024), Ny ~ U{8..64}, k ~ U[0.5, 3],
    x_t ~ U[0.3, 0.6], p0 ~ U[2, 10] bar, T0 ~ U[300, 800] K."""
    rng = np.random.default_rng(seed)
    nx = np.clip(np.rint(np.exp(rng.normal(math.log(256.0), 0.6, n))), *nx_range).astype(int)
    ny = rng.integers(ny_range[0], ny_range[1] + 1, n)
    k = rng.uniform(0.5, 3.0, n)
    xt = rng.uniform(0.3, 0.6, n)
    p0 = rng.uniform(2e5, 10e5, n)
    T0 = rng.uniform(300.0, 800.0, n)
    return [area_nozzle(int(nx[c]), int(ny[c]), float(k[c]), float(xt[c]), float(p0[c]),
                        float(T0[c])) for c in range(n)]


def closed_box(ni: int = 24, nj: int = 24, seed: int = 3, **options) -> CaseSpec:
    """A closed curvilinear box (slip walls, BC 300, on all four faces) holding a random state:
    mass and energy can only change by round-off. Options default to van Leer, RK3,
    CFL 0.4, time-accurate."""
    rng = np.random.default_rng(seed)
    x, y = np.meshgrid(np.linspace(0, 1, ni + 1), np.linspace(0, 1, nj + 1))
    x = x + 0.02 * np.sin(2 * np.pi * y)
    nodes = np.stack([x, y], axis=-1)
    prim = np.zeros((nj, ni, 4))
    prim[..., 0] = 1 + 0.1 * rng.random((nj, ni))
    prim[..., 1] = 0.1 * rng.standard_normal((nj, ni))
    prim[..., 2] = 0.1 * rng.standard_normal((nj, ni))
    prim[..., 3] = 1 + 0.1 * rng.random((nj, ni))
    blk = BlockSpec(ni, nj, nodes, prim)
    bcs = edge_records(1, ni, nj, {f: (300, {}) for f in (1, 2, 3, 4)})
    opts = dict(limiter="vanleer", n_rk=3, cfl=0.4, time_accurate=1)
    opts.update(options)
    return CaseSpec("box", [blk], bcs, opts)


def periodic_box(ni: int = 32, nj: int = 24, seed: int = 5, **options) -> CaseSpec:
    """A doubly periodic curvilinear unit square: each edge is a translational periodic seam
    (BC 201) onto the opposite edge, the grid x = X + 0.03 sin(2 pi Y), y = Y + 0.03 sin(2 pi X)
    repeats under the offsets (1, 0) and (0, 1), and the state is random. Nothing enters or
    leaves, so mass, both momenta and energy change only by round-off. Options default to
    van Leer, RK3, CFL 0.4, time-accurate."""
    rng = np.random.default_rng(seed)
    X, Y = np.meshgrid(np.linspace(0, 1, ni + 1), np.linspace(0, 1, nj + 1))
    nodes = np.stack([X + 0.03 * np.sin(2 * np.pi * Y), Y + 0.03 * np.sin(2 * np.pi * X)], axis=-1)
    prim = np.zeros((nj, ni, 4))
    prim[..., 0] = 1 + 0.1 * rng.random((nj, ni))
    prim[..., 1] = 0.2 + 0.1 * rng.standard_normal((nj, ni))
    prim[..., 2] = -0.1 + 0.1 * rng.standard_normal((nj, ni))
    prim[..., 3] = 1 + 0.1 * rng.random((nj, ni))
    blk = BlockSpec(ni, nj, nodes, prim)
    conn = dict(d11=1, d12=0, d21=0, d22=1)
    bcs = edge_records(1, ni, nj, {
        1: lambda k: (201, dict(bs=1, is_=ni, js=k, fs=2, **conn)),
        2: lambda k: (201, dict(bs=1, is_=1, js=k, fs=1, **conn)),
        3: lambda k: (201, dict(bs=1, is_=k, js=nj, fs=4, **conn)),
        4: lambda k: (201, dict(bs=1, is_=k, js=1, fs=3, **conn))})
    opts = dict(limiter="vanleer", n_rk=3, cfl=0.4, time_accurate=1)
    opts.update(options)
    return CaseSpec("periodic_box", [blk], bcs, opts)


def cell_areas(block: BlockSpec) -> np.ndarray:
    """Quadrilateral cell areas from the nodes (half the cross product of the diagonals)."""
    X, Y = block.nodes[..., 0], block.nodes[..., 1]
    d1x, d1y = X[1:, 1:] - X[:-1, :-1], Y[1:, 1:] - Y[:-1, :-1]
    d2x, d2y = X[:-1, 1:] - X[1:, :-1], Y[:-1, 1:] - Y[1:, :-1]
    return 0.5 * np.abs(d1x * d2y - d1y * d2x)


def request_case(kind: str, cells: int, rng: np.random.Generator) -> CaseSpec:
    """One served request: a planar ramp or a quasi-2D nozzle with about `cells` cells."""
    if kind == "ramp":
        nj = max(8, int(round(math.sqrt(cells / 3.0))))
        ni = max(16, int(round(cells / nj)))
        return ramp(ni, nj, seed=int(rng.integers(1 << 31)))
    nj = int(np.clip(round(math.sqrt(cells / 8.0)), 8, 256))
    ni = max(16, int(round(cells / nj)))
    return area_nozzle(ni, nj, float(rng.uniform(0.5, 3.0)), float(rng.uniform(0.3, 0.6)),
                       float(rng.uniform(2e5, 10e5)), float(rng.uniform(300.0, 800.0)))
