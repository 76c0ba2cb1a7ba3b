"""The reference's case-directory formats, for CaseSpec objects.

write_case() lays a case out the way a Q2D run directory is laid out, so that the command-line
host (q2d_b200/lib/q2d_host) or the reference binary can read it:
  input.ini            [Q2D-Parameters] / [Q2D-Physics] / [Q2D-Numerics] / [Q2D-IO] /
                       [Q2D-Sources] keys (Register_Numerics.f90:31-76,
                       Register_Sim_Param.f90:26-29, Register_IO.f90:23-39,
                       Register_Sources.f90:33, Register_Physics.f90:24)
  INPUT/bc.txt         Read_BCfile records: b, i, j, f, type, then the type's property line
                       (IO_BC.f90:163-440)
  INPUT/ic.tec         Tecplot ASCII, DATAPACKING=BLOCK, x and y nodal, rho1, u, v, p
                       cell-centred, i fastest, one zone per block (Read_IC,
                       IO_Solution.f90:38-129; test/1D/ShuOsher-LIMO3/gen_case.py:60-75)
  INPUT/block<b>_area.dat   nodal cross-section, i fastest (Lib_Source_Areavariation.f90:53-101)
  INPUT/phase.txt, INPUT/thermo.dat   one constant-cp species (the layout of test/common/Air)
read_field() reads a Tecplot BLOCK file of that layout back (the OUTPUT/field.tec the host
writes).
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

from . import _abi
from .cases import BlockSpec, CaseSpec

RUNIV = 8314.46   # docs/theory/thermo.md:56

_LIM_NAMES = {1: "minmod", 2: "vanleer", 3: "vanalbada", 4: "mc", 5: "superbee", 6: "LIMO3"}
_RIEMANN_NAMES = {0: "HLLC", 1: "HLLE", 2: "LLF", 3: "SLAU", 4: "SLAU2", 5: "HLLC+", 6: "HLLE++", 7: "HLLEM",
                  8: "HLLC Rotated", 9: "PLLF", 10: "exact", 11: "Hanel", 12: "AUSM+", 13: "AUSM+-up",
                  14: "AUSM+-up2"}
_SCHEME_NAMES = {1: "euler", 2: "RK2", 3: "RK3"}
_SOURCE_NAMES = {0: "none", 1: "axisymmetric", 2: "area_variation"}


def _fmt(x: float) -> str:
    return f"{x: .17E}"


def _ini(o: _abi.Options) -> str:
    lines = ["[Q2D-Parameters]",
             f"res-threshold = {o.res_threshold!r}",
             f"time-threshold = {o.time_threshold!r}",
             f"iter-threshold = {o.itermax}",
             "", "[Q2D-Physics]", "equations = euler",
             "", "[Q2D-Numerics]",
             f"cfl = {o.cfl!r}",
             f"cfl-rise-threshold = {o.rampa_iter}",
             f"time-scheme = {_SCHEME_NAMES[o.n_rk]}",
             f"time-accurate = {'true' if o.time_accurate else 'false'}",
             f"irs-beta = {o.irs_beta!r}",
             "integration-variables = cons"]
    if o.limiter == 0:
        lines.append("space-reconstruction = first-order")
    else:
        recon = "MUSCL-SD" if o.shock_detector else "MUSCL"
        lines += [f"space-reconstruction = {recon}", f"flux-limiter = {_LIM_NAMES[o.limiter]}"]
    if o.riemann_minf > 0.0:
        lines.append(f"riemann-options-Minf = {o.riemann_minf!r}")
    lines += [f"riemann-solver = {_RIEMANN_NAMES[o.riemann]}",
              "", "[Q2D-IO]",
              f"res-diter = {o.res_diter}",
              f"sol-diter = {o.sol_diter}",
              f"sol-dtime = {o.sol_dtime!r}",
              "", "[Q2D-Sources]",
              f"active = {_SOURCE_NAMES[o.source]}", ""]
    return "\n".join(lines)


def _dir_tok(alpha: float) -> str:
    return "normal" if alpha >= 0.5 * _abi.NORMAL_DIR else _fmt(alpha)


def _bc_lines(r: dict) -> list:
    get = lambda k, d=0.0: r.get(k, d)
    t = r["type"]
    out = [f"{r['b']:8d}{r['i']:8d}{r['j']:8d}{r['f']:8d}{t:8d}"]
    if t in (101, 201):
        vals = [r.get("bs", 0), r.get("is_", r.get("is", 0))] + [r.get(k, 0) for k in ("js", "fs", "d11", "d12", "d21", "d22")]
        out.append("".join(f"{int(v):8d}" for v in vals))
    elif t == 401:
        out.append(f"{_fmt(get('T0'))}, {_fmt(get('p0'))}, {_dir_tok(get('alpha', _abi.NORMAL_DIR))}, normal, "
                   f"{_fmt(get('rel_fac', 1.0))}, {_fmt(1.0)},")
    elif t == 405:
        out.append(f"{_fmt(get('mach'))}, {_fmt(get('T0'))}, {_fmt(get('pamb'))}, "
                   f"{_dir_tok(get('alpha', _abi.NORMAL_DIR))}, normal, {_fmt(get('rel_fac', 1.0))}, {_fmt(1.0)},")
    elif t == 406:
        out.append(f"{_fmt(get('pamb'))}, {_fmt(get('rel_fac', 1.0))},")
    return out


def write_case(cs: CaseSpec, directory, extra_ini: str = "", thermo_table=None, **option_overrides) -> Path:
    """Writes the case directory; options are the case's (make_options) with the overrides.
    extra_ini is appended to input.ini (more [Q2D-IO] keys, probe sections). thermo_table =
    (h, cp) on the knots T = 0, 1, .. K writes INPUT/thermo.dat from knot 1 on (the file's rows
    start at 1 K); without it the table holds the constant cp of gas_gamma."""
    from .solver import make_options
    o = make_options(cs, **option_overrides)
    d = Path(directory)
    (d / "INPUT").mkdir(parents=True, exist_ok=True)
    (d / "input.ini").write_text(_ini(o) + ("\n" + extra_ini if extra_ini else ""))
    with open(d / "INPUT" / "bc.txt", "w") as f:
        for r in cs.bcs:
            f.write("\n".join(_bc_lines(r)) + "\n")
    with open(d / "INPUT" / "ic.tec", "w") as f:
        f.write(' VARIABLES ="x"  "y"  "rho1"  "u"  "v"  "p"\n')
        for b, B in enumerate(cs.blocks):
            f.write(f" ZONE  T = B{b + 1}-IG, I={B.ni + 1}, J={B.nj + 1}, K=1, DATAPACKING=BLOCK, "
                    "VARLOCATION=([1-2]=NODAL,[3-6]=CELLCENTERED), SOLUTIONTIME=0.000000000000000E+000\n")
            nodes = np.asarray(B.nodes, dtype=np.float64)
            vals = [nodes[..., 0].ravel(), nodes[..., 1].ravel()]
            vals += [np.asarray(B.prim[..., v], dtype=np.float64).ravel() for v in range(4)]
            np.savetxt(f, np.concatenate(vals), fmt="% .17E")
            if B.area is not None:
                np.savetxt(d / "INPUT" / f"block{b + 1}_area.dat", np.asarray(B.area, dtype=np.float64).ravel(),
                           fmt="  %.17E")
    W = RUNIV / o.gas_R
    (d / "INPUT" / "phase.txt").write_text(f"ideal-gas phase\nair {W!r}\n")
    cp = o.gas_gamma * o.gas_R / (o.gas_gamma - 1.0)
    if thermo_table is None:
        rows = [(T, cp, cp * T) for T in (1.0, 2.0)]
    else:
        h, c = (np.asarray(t, dtype=np.float64) for t in thermo_table)
        rows = [(float(T), float(c[T]), float(h[T])) for T in range(1, len(h))]
    with open(d / "INPUT" / "thermo.dat", "w") as f:
        f.write('TITLE = "Mass Thermodynamic Properties"\n'
                'VARIABLES = "Temperature", "Cp", "Enthalpy", "Entropy", "dCp"\n'
                f'ZONE T="air"\nI={len(rows)}, F=POINT\n')
        for T, c_, h_ in rows:
            f.write(f"{T:.1f} {c_!r} {h_!r} 0.000000 0.000000\n")
    return d


def read_field(path) -> list:
    """Blocks of a Tecplot BLOCK file (x, y nodal; rho1, u, v, p cell-centred) as BlockSpec
    with nodes (nj+1, ni+1, 2) and prim (nj, ni, 4)."""
    text = Path(path).read_text().splitlines()
    blocks, k = [], 0
    while k < len(text):
        line = text[k].strip()
        k += 1
        if not line.upper().startswith("ZONE"):
            continue
        fields = {}
        for part in line[4:].replace(" ", "").split(","):
            if "=" in part:
                key, val = part.split("=", 1)
                fields[key.upper()] = val
        I, J = int(fields["I"]), int(fields["J"])
        ni, nj = I - 1, J - 1
        need = 2 * I * J + 4 * ni * nj
        vals = []
        while len(vals) < need:
            vals += [float(t.replace("D", "E").replace("d", "e")) for t in text[k].replace(",", " ").split()]
            k += 1
        a = np.array(vals)
        nn = I * J
        nodes = np.stack([a[:nn].reshape(J, I), a[nn:2 * nn].reshape(J, I)], axis=-1)
        prim = np.stack([a[2 * nn + v * ni * nj: 2 * nn + (v + 1) * ni * nj].reshape(nj, ni) for v in range(4)],
                        axis=-1)
        blocks.append(BlockSpec(ni, nj, nodes, prim))
    return blocks


def host_binary() -> Path:
    """The command-line host built next to the library (make in q2d_b200/csrc)."""
    p = _abi.LIB_DIR / "q2d_host"
    if not p.exists() or not os.access(p, os.X_OK):
        _abi.build_library(force=True)
    return p
