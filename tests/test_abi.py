"""The C ABI boundary, without a GPU: libpdot.so loads, exports every symbol
include/pdot.h declares, the ctypes mirror has the C layout, and argument
validation answers with error codes (no compute call is made)."""
import ctypes as ct
import os
import re
import subprocess

import pytest

from pdot import _abi, api, solve

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for mt in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(pdot_\w+)\s*\(", text, flags=re.M):
            names.append(mt.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "pdot_optimize" in names and "pdot_primal_pass_f64" in names


def test_library_exports_every_declared_symbol(built):
    lib = ct.CDLL(_abi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes signature table covers them all
    assert set(declared_functions()) <= set(_abi.SIGNATURES)


def test_version(built):
    assert _abi.load().pdot_version() == _abi.ABI_VERSION


STRUCTS = {
    "pdot_problem": _abi.ProblemC,
    "pdot_termination_criteria": _abi.TerminationCriteriaC,
    "pdot_restart_parameters": _abi.RestartParametersC,
    "pdot_pdhg_parameters": _abi.PdhgParametersC,
    "pdot_solver_options": _abi.SolverOptionsC,
    "pdot_solver_status": _abi.SolverStatusC,
    "pdot_convergence_information": _abi.ConvergenceInformationC,
    "pdot_iteration_stats": _abi.IterationStatsC,
    "pdot_saddle_point_output": _abi.SaddlePointOutputC,
    "pdot_batch_problem": _abi.BatchProblemC,
    "pdot_batch_output": _abi.BatchOutputC,
}


def test_ctypes_layout_matches_c(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pdot.h"', "int main(void) {"]
    expect = []
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        expect.append(ct.sizeof(cls))
        for fname, _ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append(getattr(cls, fname).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect


def test_default_parameters_match_script(built):
    lib = _abi.load()
    c = _abi.PdhgParametersC()
    lib.pdot_default_parameters(1e-4, ct.byref(c))
    p = api.marshal_params(solve.default_parameters(1e-4))
    assert bytes(c) == bytes(p)


def _problem(m=4, n=3):
    import numpy as np

    C = np.asfortranarray(np.ones((m, n)))
    return api.MarshalledProblem(api.OptimalTransportProblem(C, np.full(m, 1 / m), np.full(n, 1 / n)))


@pytest.mark.parametrize("mutate", [
    lambda p: setattr(p, "primal_importance", 0.0),
    lambda p: setattr(p, "primal_importance", float("inf")),
    lambda p: setattr(p.restart_params, "restart_frequency_if_fixed", 1),
    lambda p: setattr(p.restart_params, "artificial_restart_threshold", 0.0),
    lambda p: setattr(p.restart_params, "sufficient_reduction_for_restart", 0.95),
    lambda p: setattr(p.restart_params, "primal_weight_update_smoothing", 1.5),
    lambda p: setattr(p, "termination_evaluation_frequency", 0),
    lambda p: setattr(p, "step_size_policy", 7),
])
def test_invalid_parameters_rejected_before_any_device_work(built, mutate):
    lib = _abi.load()
    c = _abi.PdhgParametersC()
    lib.pdot_default_parameters(1e-4, ct.byref(c))
    mutate(c)
    mp = _problem()
    out = _abi.SaddlePointOutputC()
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(c), None, ct.byref(out))
    assert rc == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert _abi.last_error(lib)


def test_empty_and_null_inputs_rejected(built):
    lib = _abi.load()
    c = _abi.PdhgParametersC()
    lib.pdot_default_parameters(1e-4, ct.byref(c))
    out = _abi.SaddlePointOutputC()
    mp = _problem()
    empty = _abi.ProblemC(0, 3, mp.c.cost_matrix, mp.c.source_distribution, mp.c.target_distribution)
    assert lib.pdot_optimize(ct.byref(empty), ct.byref(c), None, ct.byref(out)) == _abi.PDOT_ERR_INVALID_ARGUMENT
    nullc = _abi.ProblemC(4, 3, None, mp.c.source_distribution, mp.c.target_distribution)
    assert lib.pdot_optimize(ct.byref(nullc), ct.byref(c), None, ct.byref(out)) == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert lib.pdot_optimize(ct.byref(mp.c), ct.byref(c), None, None) == _abi.PDOT_ERR_INVALID_ARGUMENT


def test_no_device_is_an_error_code_not_a_crash(built):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = _abi.load()
    c = _abi.PdhgParametersC()
    lib.pdot_default_parameters(1e-4, ct.byref(c))
    mp = _problem()
    out = _abi.SaddlePointOutputC()
    assert lib.pdot_optimize(ct.byref(mp.c), ct.byref(c), None, ct.byref(out)) == _abi.PDOT_ERR_NO_DEVICE
    with pytest.raises(_abi.PdotError):
        api.optimize(solve.default_parameters(1e-4), api.OptimalTransportProblem(
            mp.C, mp.a, mp.b))


def test_python_validation_mirrors_reference():
    with pytest.raises(AssertionError):
        api.construct_restart_parameters(api.ADAPTIVE_KKT, api.KKT_GREEDY, 1, 0.36, 0.1, 0.9, 0.5)
    with pytest.raises(AssertionError):
        api.construct_restart_parameters(api.ADAPTIVE_KKT, api.KKT_GREEDY, 1000, 0.36, 0.5, 0.4, 0.5)
    params = solve.default_parameters(1e-4)
    params.primal_importance = -1.0
    with pytest.raises(ValueError):
        api.optimize(params, api.OptimalTransportProblem(*_problem_arrays()))


def _problem_arrays():
    import numpy as np

    return np.ones((2, 2)), np.full(2, 0.5), np.full(2, 0.5)
