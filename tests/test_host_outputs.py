"""Solution outputs and probes of the command-line host (q2d_host).

* Probes ([Q2D-Probes] probe<n> = name, a section per probe; IO_Probes.f90, Register_IO.f90:
  44-82): parsed with their variables, frequencies and cell, placed at the nearest grid node when
  given by position; on the GPU, the reference's prandtl-meyer case (test/2D/euler/prandtl-meyer)
  written with its probe 'exit' (Mach every 100 iterations at cell 1 50 33) reaches the exit
  Mach number of its check.py, the Prandtl-Meyer expansion of Mach 2 by 34.971 degrees, within
  the case's 0.5 %.
* Write_Solution (Wrap_Postprocess.f90:104-125, IO_Solution.f90:234-326): sol-overwrite = false
  numbers the intermediate solutions field1, field2, ...; sol-format = vtk ascii / vtk raw writes
  VTK XML structured grids (OUTPUT/vtk/<stem>_Block<b>.vts, index OUTPUT/<stem>.vtm) holding the
  same values as the Tecplot output.
"""
import json
import re
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from q2d_b200 import cases, refio
from tests.helpers import prandtl_meyer_case, prandtl_meyer_exit_mach


def host(*args, check=True):
    r = subprocess.run([str(refio.host_binary()), *map(str, args)], capture_output=True, text=True, timeout=900)
    if check and r.returncode != 0:
        raise AssertionError(f"q2d_host {args}: rc={r.returncode}\n{r.stdout}\n{r.stderr}")
    return r


PROBES = """[Q2D-Probes]
probe1 = exit
probe2 = corner

[exit]
variables = M
diter = 100
index-position = 1 50 33

[corner]
variables = rho(1) u v p T M
diter = 250
position = 0.5 0.02
"""


def test_probes_parsed_and_placed(tmp_path):
    cs = prandtl_meyer_case()
    refio.write_case(cs, tmp_path, extra_ini=PROBES)
    info = json.loads(host(tmp_path, "--check").stdout)
    exit_p, corner = info["probes"]
    assert exit_p == {"file": "exit", "variables": ["M"], "diter": 100, "dtime": 1e30, "cell": [1, 50, 33]}
    assert corner["variables"] == ["rho(1)", "u", "v", "p", "T", "M"] and corner["diter"] == 250
    # nearest node (i = 1..ni, j = 0..nj) to the position, as Place does
    nodes = cs.blocks[0].nodes
    d = np.hypot(nodes[:, 1:, 0] - 0.5, nodes[:, 1:, 1] - 0.02)
    j, i = np.unravel_index(np.argmin(d), d.shape)
    assert corner["cell"] == [1, int(i) + 1, max(int(j), 1)]
    assert info["sol_format"] == "tecplot ascii" and info["sol_overwrite"] == 1


def test_solution_format_keys(tmp_path):
    cs = cases.ramp(20, 6, seed=3)
    refio.write_case(cs, tmp_path, extra_ini="[Q2D-IO]\nsol-format = vtk raw\nsol-overwrite = false\n")
    info = json.loads(host(tmp_path, "--check").stdout)
    assert info["sol_format"] == "vtk raw" and info["sol_overwrite"] == 0 and not info["unsupported"]
    refio.write_case(cs, tmp_path, extra_ini="[Q2D-IO]\nsol-format = tecplot binary\n")
    info = json.loads(host(tmp_path, "--check").stdout)
    assert info["unsupported"] == ["[Q2D-IO] sol-format = tecplot binary"]


@pytest.mark.gpu
def test_prandtl_meyer_exit_probe(tmp_path):
    cs = prandtl_meyer_case()
    refio.write_case(cs, tmp_path, extra_ini=PROBES)
    host(tmp_path, "--steps-per-call", 500, "--quiet")
    hist = np.loadtxt(tmp_path / "OUTPUT" / "residuals.dat")
    last = int(hist[-1, 0])   # the run ends on res-threshold or at iter-threshold
    lines = [ln.split() for ln in (tmp_path / "OUTPUT" / "exit.txt").read_text().splitlines() if ln.strip()]
    iters = [int(t[0]) for t in lines]
    # every 100 iterations, but not on the last one (TODO = 3 writes the solution, not the probes)
    assert iters == list(range(100, last, 100)) and iters, (iters, last)
    mach = float(lines[-1][1])
    m2 = prandtl_meyer_exit_mach()
    assert abs(mach - m2) / m2 <= 0.005, (mach, m2)
    corner = [ln.split() for ln in (tmp_path / "OUTPUT" / "corner.txt").read_text().splitlines() if ln.strip()]
    assert [int(t[0]) for t in corner] == list(range(250, last, 250)) and all(len(t) == 7 for t in corner)
    field = refio.read_field(tmp_path / "OUTPUT" / "field.tec")[0].prim
    assert np.all(field[..., 0] > 0) and np.all(field[..., 3] > 0)


def _read_vts(path):
    raw = path.read_bytes()
    head, _, tail = raw.partition(b"<AppendedData")
    text = head.decode() + ("</VTKFile>" if tail else "")   # the XML part before the raw block
    root = ET.fromstring(text if tail else raw.decode())
    blob = tail[tail.index(b"_") + 1:] if tail else b""
    out = {}
    for da in root.iter("DataArray"):
        name = da.get("Name") or "Points"
        if da.get("format") == "appended":
            off = int(da.get("offset"))
            n = int(np.frombuffer(blob[off:off + 8], dtype="<u8")[0])
            out[name] = np.frombuffer(blob[off + 8:off + 8 + n], dtype="<f8")
        else:
            out[name] = np.array([float(x) for x in da.text.split()])
    return root, out


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["vtk ascii", "vtk raw"])
def test_numbered_and_vtk_solutions(tmp_path, fmt):
    cs = cases.ramp(40, 12, seed=5)
    tec = tmp_path / "tec"
    vtk = tmp_path / "vtk"
    refio.write_case(cs, tec, itermax=30, sol_diter=10, extra_ini="[Q2D-IO]\nsol-overwrite = false\n")
    refio.write_case(cs, vtk, itermax=30, sol_diter=10,
                     extra_ini=f"[Q2D-IO]\nsol-overwrite = false\nsol-format = {fmt}\n")
    host(tec, "--quiet", "--steps-per-call", 7)
    host(vtk, "--quiet", "--steps-per-call", 7)
    names = sorted(p.name for p in (tec / "OUTPUT").glob("field*.tec"))
    assert names == ["field.tec", "field1.tec", "field2.tec"]   # IO at 10, 20; the end at 30
    stems = sorted(p.stem for p in (vtk / "OUTPUT").glob("field*.vtm"))
    assert stems == ["field", "field1", "field2"]
    for stem in stems:
        t = refio.read_field(tec / "OUTPUT" / f"{stem}.tec")[0]
        vtm = ET.parse(vtk / "OUTPUT" / f"{stem}.vtm").getroot()
        files = [d.get("file") for d in vtm.iter("DataSet")]
        assert files == [f"vtk/{stem}_Block1.vts"]
        root, arr = _read_vts(vtk / "OUTPUT" / files[0])
        ext = root.find("StructuredGrid").get("WholeExtent").split()
        assert [int(x) for x in ext] == [0, cs.blocks[0].ni, 0, cs.blocks[0].nj, 0, 0]
        pts = arr["Points"].reshape(-1, 3)
        assert np.array_equal(pts[:, :2].reshape(t.nodes.shape), t.nodes)
        for k, name in enumerate(["rho(1)", "u", "v", "p"]):
            assert np.array_equal(arr[name].reshape(t.prim.shape[:2]), t.prim[..., k]), (stem, name)
        T = arr["T"].reshape(t.prim.shape[:2])
        np.testing.assert_allclose(T, t.prim[..., 3] / (t.prim[..., 0] * 287.0), rtol=1e-14)
        assert re.search(r"TIME", (vtk / "OUTPUT" / files[0]).read_bytes()[:2000].decode(errors="ignore"))
