"""The files of scripts/solve.jl:91-120 as the reference writes them: vectors
one Float64 per line in Julia's text form, and the solve logs as JSON3
writes a SolveLog (compact, fields in declaration order, enums by name,
floats in Julia's shortest form)."""
import gzip
import json
import math
import os

import numpy as np
import pytest

import pdot
from pdot import api, instances, solve


@pytest.mark.parametrize("x,text", [
    (0.25, "0.25"), (0.1, "0.1"), (3.0, "3.0"), (-2.0, "-2.0"), (0.0, "0.0"), (-0.0, "-0.0"),
    (0.0001, "0.0001"), (1e-5, "1.0e-5"), (1.5e-7, "1.5e-7"), (5e-324, "5.0e-324"),
    (100000.0, "100000.0"), (999999.0, "999999.0"), (1e6, "1.0e6"), (1234567.0, "1.234567e6"),
    (123456789.0, "1.23456789e8"), (1e22, "1.0e22"), (12.5, "12.5"), (0.001234, "0.001234"),
    (math.inf, "Inf"), (-math.inf, "-Inf"), (math.nan, "NaN"),
])
def test_julia_float_text(x, text):
    assert solve.julia_float_str(x) == text
    if math.isfinite(x):
        assert float(text) == x  # shortest round-trip digits


def test_solve_log_json_is_compact_json3_text():
    log = api.SolveLog()
    log.instance_name = "c1"
    log.iteration_count = 640
    log.solve_time_sec = 1e-5
    log.solution_type = api.PointType.POINT_TYPE_AVERAGE_ITERATE
    text = solve.solve_log_json(log)
    assert text.startswith('{"instance_name":"c1","command_line_invocation":"",'
                           '"termination_reason":"TERMINATION_REASON_UNSPECIFIED","termination_string":"",'
                           '"iteration_count":640,"solve_time_sec":1.0e-5,"solution_stats":{')
    assert ", " not in text and '": ' not in text
    assert '"solution_type":"POINT_TYPE_AVERAGE_ITERATE","iteration_stats":[]}' in text
    parsed = json.loads(text)
    assert parsed["solve_time_sec"] == 1e-5


def test_vector_file_is_column_major_julia_text(tmp_path):
    X = np.asfortranarray([[1.0, 2.5e-6], [3e6, -0.5]])
    f = tmp_path / "v.txt"
    solve.write_vector_to_file(str(f), X)
    assert f.read_text() == "1.0\n3.0e6\n2.5e-6\n-0.5\n"


def _julia_json(text):
    """json.loads of JSON3 text with allow_inf (bare Inf / -Inf / NaN)."""
    import re

    text = re.sub(r'(?<=[:\[,])(-?)Inf(?=[,\]}])', r'\1Infinity', text)
    return json.loads(text)


def test_julia_json_reader_reads_non_finite_values():
    log = api.SolveLog()
    log.solve_time_sec = math.inf
    text = solve.solve_log_json(log)
    assert '"solve_time_sec":Inf,' in text
    assert _julia_json(text)["solve_time_sec"] == math.inf


@pytest.mark.gpu
def test_solve_instance_and_output_writes_the_scripts_files(cuda, tmp_path):
    prob = instances.uniform_sqeuclid(30, 20, seed=1)
    out = pdot.solve_instance_and_output(str(tmp_path), "t", prob, tolerance=1e-4)
    names = sorted(os.listdir(tmp_path))
    assert names == ["t_dual.txt", "t_full_log.json.gz", "t_primal.txt", "t_primal_rounded.txt", "t_summary.json"]
    summary = _julia_json((tmp_path / "t_summary.json").read_text())
    assert summary["termination_reason"] == "TERMINATION_REASON_OPTIMAL"
    assert summary["iteration_count"] == out.iteration_count and summary["iteration_stats"] == []
    with gzip.open(tmp_path / "t_full_log.json.gz", "rt") as io:
        full = _julia_json(io.read())
    assert len(full["iteration_stats"]) == len(out.iteration_stats)
    primal = np.loadtxt(tmp_path / "t_primal.txt")
    np.testing.assert_array_equal(primal, out.primal_solution.ravel(order="F"))
    dual = np.loadtxt(tmp_path / "t_dual.txt")
    assert dual.size == 50
