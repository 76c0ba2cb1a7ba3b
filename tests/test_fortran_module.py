"""The shipped Fortran interface module (include/q2d_gpu_m.f90) against the C header: no Fortran
compiler exists here, so its text is parsed. Every bind(c) derived type must list the fields of
its C struct in the same order with the same kinds (checked as ctypes layouts: offsets and
size), and the module must declare an interface for every entry point of include/q2d_gpu.h."""
import ctypes as C
import re
from pathlib import Path

from q2d_b200 import _abi
from tests.test_abi import declared_functions

MOD = Path(__file__).resolve().parents[1] / "include" / "q2d_gpu_m.f90"
KINDS = {"integer(c_int)": C.c_int, "integer(c_long_long)": C.c_longlong, "real(c_double)": C.c_double,
         "real(c_float)": C.c_float}


def module_text():
    return "\n".join(line.split("!")[0] for line in MOD.read_text().splitlines())


def bind_c_types():
    txt = module_text()
    out = {}
    for name, body in re.findall(r"type\s*,\s*bind\(c\)\s*::\s*(\w+)(.*?)end\s+type", txt, flags=re.S | re.I):
        fields = []
        for line in body.splitlines():
            if "::" not in line:
                continue
            kind, names = (x.strip() for x in line.split("::", 1))
            ctype = KINDS[kind.lower().replace(" ", "")]
            for item in re.split(r",\s*(?![^()]*\))", names):
                m = re.fullmatch(r"(\w+)\s*(?:\((\d+)\))?", item.strip())
                nm, cnt = m.group(1), int(m.group(2) or 1)
                fields.append((nm.lower(), ctype * cnt if cnt > 1 else ctype))
        out[name.lower()] = fields
    return out


def layout(fields):
    S = type("S", (C.Structure,), {"_fields_": fields})
    return C.sizeof(S), [(n, getattr(S, n).offset, getattr(S, n).size) for n, _ in fields]


def test_derived_types_match_the_c_structs():
    types = bind_c_types()
    pairs = {"q2d_options": _abi.Options, "q2d_bc_rec": _abi.BCRec, "q2d_step_info": _abi.StepInfo}
    assert set(pairs) <= set(types)
    for fname, cls in pairs.items():
        ref = [(("is" if n == "is_" else n).lower(), t) for n, t in cls._fields_]
        got = types[fname]
        assert [n for n, _ in got] == [n for n, _ in ref], fname
        assert layout(got) == layout(ref), fname


def test_module_declares_every_entry_point():
    txt = module_text()
    declared = set(re.findall(r"(?:function|subroutine)\s+(q2d_\w+)\s*\(", txt, flags=re.I))
    assert declared == set(declared_functions())


def test_module_constants_match_the_header():
    hdr = (Path(__file__).resolve().parents[1] / "include" / "q2d_gpu.h").read_text()
    cdefs = dict(re.findall(r"#define\s+(Q2D_\w+)\s+(\d+)", hdr))
    fdefs = dict(re.findall(r"(Q2D_\w+)\s*=\s*(\d+)", module_text()))
    assert fdefs, "no constants parsed"
    for k, v in fdefs.items():
        assert cdefs.get(k) == v, k
