"""The exec command line (opengpop_b200/bin/gpop_exec): the reference's JSON contract
(exec/main.cpp:28-107). CPU tests cover argument handling and JSON parsing; GPU tests compare the
CLI's output with the library call it wraps."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "opengpop_b200", "bin", "gpop_exec")

START = {"Year": 2023, "Month": 4, "Day": 29, "Hour": 22, "Min": 59, "Sec": 42.0}


def _run(*args, cwd=None):
    return subprocess.run([EXE, *args], capture_output=True, text=True, cwd=cwd, timeout=600)


def test_cli_requires_subcommand_and_input():
    assert _run().returncode == 109
    assert _run("orbit").returncode == 109
    assert _run("propagate").returncode == 109
    r = _run("propagate", "-i", "/nonexistent.json")
    assert r.returncode == 105 and "does not exist" in r.stderr


def test_cli_rejects_malformed_json(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{"propagationStart": {"Year": 2023,, }')
    r = _run("propagate", "-i", str(p))
    assert r.returncode == 1 and "JSON parse error" in r.stderr
    p.write_text(json.dumps({"propagationSeconds": 60, "positions": [], "velocities": []}))
    r = _run("propagate", "-i", str(p))
    assert r.returncode == 1 and "propagationStart" in r.stderr


def _write_input(tmp_path, r, v, seconds, sets=None):
    d = {"propagationStart": START, "propagationSeconds": seconds,
         "positions": np.asarray(r).tolist(), "velocities": np.asarray(v).tolist()}
    if sets is not None:
        d["setIndices"] = [int(s) for s in sets]
    p = tmp_path / "in.json"
    p.write_text(json.dumps(d))
    return p


@pytest.mark.gpu
def test_cli_propagate_matches_library(tmp_path):
    import opengpop_b200 as G
    # the reference's sample input: two 6878 km orbits (data/sat_data.json layout)
    r0 = np.array([[6878136.3, 0.0, 0.0], [-6878136.3, 0.0, 0.0]])
    v0 = np.array([[0.0, 7612.6081732238688, 0.0], [0.0, -10040.175, 0.0]])
    inp = _write_input(tmp_path, r0, v0, 46800)
    out = tmp_path / "out.json"
    r = _run("propagate", "-i", str(inp), "-o", str(out))
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    d = json.loads(text)
    assert sorted(d) == ["positionsEnd", "positionsStart", "propagationSeconds",
                         "propagationStart", "velocitiesEnd", "velocitiesStart"]
    assert text.startswith('{\n    "positionsEnd": [\n        [\n')
    ctx = G.Context()
    re, ve = ctx.propagate((2023, 4, 29, 22, 59, 42.0), 46800 / 1560, 1560, r0, v0)
    assert np.array_equal(np.array(d["positionsEnd"]), re)
    assert np.array_equal(np.array(d["velocitiesEnd"]), ve)
    assert d["propagationStart"] == START and d["propagationSeconds"] == 46800


@pytest.mark.gpu
def test_cli_closest_approach_matches_library(tmp_path):
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(12, seed=31)
    r0[8:12] = r0[0:4] + np.array([700.0, 300.0, -100.0])
    v0[8:12] = v0[0:4]
    sets = [0] * 6 + [1] * 6
    inp = _write_input(tmp_path, r0, v0, 3600, sets)
    out = tmp_path / "ca.json"
    r = _run("closest-approach", "-i", str(inp), "-o", str(out))
    assert r.returncode == 0, r.stderr
    d = json.loads(out.read_text())
    recs = d["closestApproaches"]
    assert len(recs) == 36
    assert sorted(recs[0]) == ["distance", "objectIndex1", "objectIndex2", "positionAx",
                               "positionAy", "positionAz", "positionBx", "positionBy",
                               "positionBz", "time"]
    ctx = G.Context()
    ca = ctx.closest_approach((2023, 4, 29, 22, 59, 42.0), 30.0, r0, v0, sets)
    ca.propagate(120)
    lib = ca.find()
    assert [(x["objectIndex1"], x["objectIndex2"]) for x in recs] == \
        [(x.object_index1, x.object_index2) for x in lib]
    assert np.array_equal([x["distance"] for x in recs], [x.distance for x in lib])
    # --threshold keeps the pairs below it
    r = _run("closest-approach", "-i", str(inp), "-o", str(out), "--threshold", "5000")
    assert r.returncode == 0
    d = json.loads(out.read_text())
    assert all(x["distance"] < 5000 for x in d["closestApproaches"])
    assert len(d["closestApproaches"]) == sum(1 for x in lib if x.distance < 5000)


def test_streaming_json_writer_matches_whole_document(tmp_path):
    # the closest-approach output is written record by record; the bytes must equal those of the
    # whole-document writer (the reference's dump(4) layout)
    import subprocess
    exe = str(tmp_path / "json_stream_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "opengpop_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "json_stream_check.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    assert subprocess.run([exe]).returncode == 0


def _nlohmann_include():
    """Directory holding nlohmann/json.hpp 3.11.3 in this Python environment (a vendored copy in
    cudnn_frontend's package), or None."""
    import glob
    import site
    import sysconfig
    roots = set(site.getsitepackages() + [sysconfig.get_paths()["purelib"]])
    for root in sorted(roots):
        for hdr in glob.glob(os.path.join(root, "**", "nlohmann", "json.hpp"), recursive=True):
            with open(hdr, errors="replace") as f:
                head = f.read(4000)
            if "NLOHMANN_JSON_VERSION_MINOR 11" in head and "NLOHMANN_JSON_VERSION_PATCH 3" in head:
                return os.path.dirname(os.path.dirname(hdr))
    return None


def test_json_writer_bytes_equal_nlohmann(tmp_path):
    # The reference writes its output with nlohmann::json's dump(4) (exec/main.cpp:87-88,100-101).
    # The CLI's writer must give the same bytes: numbers (edge values and ~1.4 million random
    # doubles), string escapes, and whole propagate / closest-approach documents, streamed or not.
    import subprocess
    inc = _nlohmann_include()
    if inc is None:
        pytest.skip("nlohmann/json 3.11.3 header not found in this environment")
    exe = str(tmp_path / "json_nlohmann_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "opengpop_b200", "csrc"),
                    "-I", inc, os.path.join(ROOT, "tests", "cpp", "json_nlohmann_check.cpp"), "-o",
                    exe], check=True, capture_output=True, text=True)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and p.stdout.strip().endswith("ok"), p.stdout[-3000:]


def test_json_writer_power_table():
    # the writer's cached powers of ten: 10^k (k = -300, -292, ..., 324) rounded to nearest as a
    # 64-bit significand with its top bit set, times 2^e; recomputed here with exact rationals
    import re
    from fractions import Fraction
    text = open(os.path.join(ROOT, "opengpop_b200", "csrc", "json.h")).read()
    rows = re.findall(r"\{ 0x([0-9A-F]{16})ULL, (-?\d+), (-?\d+) \}", text)
    assert [int(k) for _, _, k in rows] == list(range(-300, 325, 8))
    for f_hex, e, k in rows:
        f, e, k = int(f_hex, 16), int(e), int(k)
        assert 2 ** 63 <= f < 2 ** 64
        exact = Fraction(10) ** k / Fraction(2) ** e
        assert abs(exact - f) <= Fraction(1, 2), k
