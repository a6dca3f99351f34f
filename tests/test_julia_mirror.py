"""The Julia module's C mirrors (pdot.jl_b200/julia/PDOT.jl) against the C ABI.

No Julia toolchain runs here, so the Julia struct definitions are read as text:
each field's C size and alignment follow from its Julia type (isbits structs
have the C layout), and the resulting offsets and sizes must equal those of
the ctypes mirrors, which tests/test_abi.py checks against the compiled
header. The Julia function bodies are not exercised."""
import ctypes as ct
import os
import re

import pytest

from pdot import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "pdot.jl_b200", "julia", "PDOT.jl")

PRIM = {"Int32": (4, 4), "Int64": (8, 8), "Float64": (8, 8), "Float32": (4, 4), "Cint": (4, 4)}


def julia_structs():
    text = open(JL).read()
    out = {}
    for mt in re.finditer(r"^(?:mutable )?struct (C[A-Z]\w*)[ \t]*(?:#[^\n]*)?\n(.*?)^end", text, flags=re.M | re.S):
        fields = []
        for line in mt.group(2).splitlines():
            line = line.split("#")[0].strip()
            fm = re.match(r"(\w+)::(.+)$", line)
            if fm:
                fields.append((fm.group(1), fm.group(2).strip()))
        out[mt.group(1)] = fields
    return out


def layout(tname, structs):
    """(size, align, {field: offset}) of a Julia type in C layout."""
    if tname in PRIM:
        return PRIM[tname][0], PRIM[tname][1], {}
    if tname.startswith("Ptr{"):
        return 8, 8, {}
    m = re.match(r"NTuple\{(\d+),\s*(\w+)\}", tname)
    if m:
        s, a, _ = layout(m.group(2), structs)
        return s * int(m.group(1)), a, {}
    fields = structs[tname]
    off, align, offs = 0, 1, {}
    for name, ft in fields:
        s, a, _ = layout(ft, structs)
        off = (off + a - 1) // a * a
        offs[name] = off
        off += s
        align = max(align, a)
    return (off + align - 1) // align * align, align, offs


MIRRORS = {
    "CProblem": _abi.ProblemC,
    "CTerminationCriteria": _abi.TerminationCriteriaC,
    "CRestartParameters": _abi.RestartParametersC,
    "CPdhgParameters": _abi.PdhgParametersC,
    "CConvergenceInformation": _abi.ConvergenceInformationC,
    "CIterationStats": _abi.IterationStatsC,
    "COutput": _abi.SaddlePointOutputC,
    "CSolverOptions": _abi.SolverOptionsC,
    "CBatchProblem": _abi.BatchProblemC,
    "CBatchOutput": _abi.BatchOutputC,
}


def test_every_julia_mirror_is_checked():
    assert set(julia_structs()) == set(MIRRORS)


@pytest.mark.parametrize("jname", sorted(MIRRORS))
def test_julia_mirror_layout_matches_c(jname):
    structs = julia_structs()
    cls = MIRRORS[jname]
    size, _, offs = layout(jname, structs)
    assert size == ct.sizeof(cls), (jname, size, ct.sizeof(cls))
    cfields = {name for name, _ in cls._fields_}
    checked = 0
    for name, off in offs.items():
        if name in cfields:
            assert off == getattr(cls, name).offset, (jname, name)
            checked += 1
    if jname == "CConvergenceInformation":  # 16 doubles gathered in one NTuple
        assert offs["values"] == getattr(cls, cls._fields_[1][0]).offset
    else:
        assert checked == len(cls._fields_), (jname, cfields - set(offs))
