"""Generates the committed golden fixtures of tests/golden from the reference tree.

Run in a container that has the reference checkout (it is not needed afterwards):
    python tests/golden/make_golden.py /path/to/open-hydra-Q2D

Fixtures written (all small text/npz files):
  shuosher_<lim>.txt  outputs of the reference binary for the Shu-Osher problem at N=400,
                      t=1.8, HLLC, RK3, CFL 0.5, one per limiter (copied verbatim from
                      test/1D/ShuOsher-LIMO3/reference/baseline_{iord,minmod,vanleer,mc}.dat)
  sod79_exact.txt     exact Sod solution at t=0.2 (test/1D/Sod79/reference/exact.txt)
  riemann_exact.npz   exact Riemann solutions sampled at cell centres for the seeded 1-D
                      Riemann workloads, from the reference's own exact solver
                      (test/common/pycheck/q2d_exact1d.py:riemann_exact, imported, not copied)
  chang_nozzle.npz    the reference's chang-nozzle case (test/2D/euler/chang-nozzle): its grid
                      nodes and initial state read from INPUT/ic.tec, the stagnation values of
                      its BC 401 records (INPUT/bc.txt), and Chang's (1996) Mach number along the
                      axis and the wall that its check.py compares against (reference/ref1.dat,
                      ref2.dat)
  prandtl_meyer.npz   the reference's prandtl-meyer case (test/2D/euler/prandtl-meyer): its grid,
                      initial state and bc.txt records (type; M, T, p of the supersonic inflow)
  ramp_channel.npz    the reference's ramp-channel case (test/2D/euler/ramp-channel): its grid
                      nodes and initial state read from INPUT/ic.tec and the Mach number,
                      temperature and pressure of its BC 405 records (INPUT/bc.txt)
  planar_nozzle_residuals.txt   iteration and density residual of every line the reference
                      binary printed while solving its planar-nozzle case (IRS beta 0.5,
                      stagnation inflow, area-variation source; test/2D/euler/planar-nozzle/
                      solve.log), the last line being the iteration that met res-threshold
"""
import importlib.util
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    for lim in ("iord", "minmod", "vanleer", "mc"):
        shutil.copyfile(ref / f"test/1D/ShuOsher-LIMO3/reference/baseline_{lim}.dat",
                        HERE / f"shuosher_{lim}.txt")
    shutil.copyfile(ref / "test/1D/Sod79/reference/exact.txt", HERE / "sod79_exact.txt")

    spec = importlib.util.spec_from_file_location(
        "q2d_exact1d", ref / "test/common/pycheck/q2d_exact1d.py")
    ex = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ex)
    from q2d_b200 import cases

    out = {}
    for tag, seed, ni in (("cfg1", cases.BASE_SEED, 1024), ("s1", 11, 256), ("s2", 12, 256)):
        cs = cases.riemann_1d(ni=ni, seed=seed)
        rl, ul, pl, rr, ur, pr = cs.meta["states"]
        xc = 0.5 * (np.linspace(0, 1, ni + 1)[:-1] + np.linspace(0, 1, ni + 1)[1:])
        sol = ex.riemann_exact(xc, cs.meta["t_end"], 0.5, rl, ul, pl, rr, ur, pr, 1.4)
        rho, u, p = sol["rho"], sol["u"], sol["p"]
        out[f"{tag}_states"] = np.array([rl, ul, pl, rr, ur, pr, ni, seed, cs.meta["t_end"]])
        out[f"{tag}_rho"], out[f"{tag}_u"], out[f"{tag}_p"] = rho, u, p
    # Toro test 1 (Sod) known answer of the exact solver: p* = 0.30313, u* = 0.92745
    sol = ex.riemann_exact(np.array([0.5]), 0.2, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4)
    out["toro1_pstar_ustar"] = np.array([sol["pstar"], sol["ustar"]])
    np.savez(HERE / "riemann_exact.npz", **out)
    from q2d_b200 import refio
    cdir = ref / "test/2D/euler/chang-nozzle"
    blk = refio.read_field(cdir / "INPUT" / "ic.tec")[0]
    props = None
    lines = (cdir / "INPUT" / "bc.txt").read_text().splitlines()
    for k, line in enumerate(lines):
        t = line.split()
        if len(t) == 5 and t[4] == "401":
            vals = lines[k + 1].replace(",", " ").split()
            cur = (float(vals[0]), float(vals[1]))
            assert props is None or props == cur
            props = cur
    np.savez_compressed(HERE / "chang_nozzle.npz", nodes=blk.nodes, prim=blk.prim, T0_p0=np.array(props),
                        axis_mach=np.loadtxt(cdir / "reference" / "ref1.dat"),
                        wall_mach=np.loadtxt(cdir / "reference" / "ref2.dat"))
    rdir = ref / "test/2D/euler/ramp-channel"
    blk = refio.read_field(rdir / "INPUT" / "ic.tec")[0]
    props = None
    lines = (rdir / "INPUT" / "bc.txt").read_text().splitlines()
    for k, line in enumerate(lines):
        t = line.split()
        if len(t) == 5 and t[4] == "405":
            vals = lines[k + 1].replace(",", " ").split()
            cur = (float(vals[0]), float(vals[1]), float(vals[2]))
            assert props is None or props == cur
            props = cur
    np.savez_compressed(HERE / "ramp_channel.npz", nodes=blk.nodes, prim=blk.prim, mach_T_p=np.array(props))
    pdir = ref / "test/2D/euler/prandtl-meyer"
    blk = refio.read_field(pdir / "INPUT" / "ic.tec")[0]
    recs = []
    lines = (pdir / "INPUT" / "bc.txt").read_text().splitlines()
    for k, line in enumerate(lines):
        t = line.split()
        if len(t) == 5:
            b, i, j, f, typ = (int(x) for x in t)
            props = (0.0, 0.0, 0.0)
            if typ == 405:
                vals = lines[k + 1].replace(",", " ").split()
                props = (float(vals[0]), float(vals[1]), float(vals[2]))
            recs.append((b, i, j, f, typ) + props)
    np.savez_compressed(HERE / "prandtl_meyer.npz", nodes=blk.nodes, prim=blk.prim, bcs=np.array(recs))
    rows = []
    for line in (ref / "test/2D/euler/planar-nozzle/solve.log").read_text().splitlines():
        if "| Iter =" in line and "Density residual" in line:
            it = int(line.split("Iter =")[1].split("|")[0])
            res = float(line.split("Density residual =")[1].replace("D", "E"))
            rows.append((it, res))
    np.savetxt(HERE / "planar_nozzle_residuals.txt", np.array(rows), fmt=["%d", "%.6E"],
               header="iteration density_residual (reference binary, test/2D/euler/planar-nozzle/solve.log)")
    print("written:", sorted(p.name for p in HERE.iterdir() if p.suffix in (".txt", ".npz")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
