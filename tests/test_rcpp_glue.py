"""The Rcpp glue a maintainer adds to rwig (rwig_b200/rcpp/rwig_b200_glue.cpp)
compiled outside R against a stand-in Rcpp.h (tests/rcpp_stub/), linked to the
engine and run: on a machine without a GPU every GPU branch must turn the
engine's error into an R error (Rcpp::stop); on a GPU its results must equal
the Python API's on the same inputs."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "rwig_b200")


def _build(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIB_DIR, "librwig_b200.so")):
        pytest.skip("engine library not built")
    exe = str(tmp_path / "glue_main")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "tests", "rcpp_stub"),
                    "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "rcpp_stub", "glue_main.cpp"),
                    os.path.join(ROOT, "rwig_b200", "rcpp", "rwig_b200_glue.cpp"),
                    "-L", LIB_DIR, "-lrwig_b200", f"-Wl,-rpath,{LIB_DIR}"], check=True)
    return exe


def _run(exe):
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.strip().splitlines()
    assert [ln.split()[1] for ln in out] == ["sinkhorn_vanilla", "sinkhorn_log", "barycenter_parallel",
                                            "barycenter_log", "wdl"], out
    return out


def test_glue_compiles_links_and_raises_r_errors_without_a_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the gpu test below covers the call path")
    for line in _run(_build(tmp_path)):
        assert line.startswith("error ") and "device" in line, line


def _inputs():
    n, S = 24, 3
    i = np.arange(n)
    a = (1.0 + i % 5) / (3.0 * n)
    b = (1.0 + i % 7) / (4.0 * n)
    C = ((i[:, None] - i[None, :]) / 24.0) ** 2
    s = np.arange(S)
    A = (1.0 + (i[:, None] + s[None, :]) % 4) / (2.5 * n)
    w = np.full(S, 1.0 / 3)
    be = np.full(n, 1.0 / n)
    return a, b, C, A, w, be


@pytest.mark.gpu
def test_glue_results_equal_the_python_api(tmp_path):
    import rwig_b200 as rw
    lines = {ln.split()[1]: ln.split() for ln in _run(_build(tmp_path))}
    assert all(v[0] == "ok" for v in lines.values()), lines
    a, b, C, A, w, be = _inputs()
    r = rw.sinkhorn(a, b, C, {"reg": 0.1, "method": "vanilla", "with_grad": True, "max_iter": 1000,
                              "zero_tol": 1e-9})
    assert int(lines["sinkhorn_vanilla"][2]) == r["return_status"] and float(lines["sinkhorn_vanilla"][4]) == r["loss"]
    r = rw.sinkhorn(a, b, C, {"reg": 0.05, "method": "log", "max_iter": 1000, "zero_tol": 1e-9})
    assert int(lines["sinkhorn_log"][3]) == r["iter"] and float(lines["sinkhorn_log"][4]) == r["loss"]
    for method in ("parallel", "log"):
        r = rw.barycenter(A, C, w, be, {"reg": 0.1, "method": method, "with_grad": True, "max_iter": 20,
                                        "zero_tol": 0.0})
        ln = lines[f"barycenter_{method}"]
        assert int(ln[2]) == r["return_status"] == 1 and int(ln[3]) == 20 and float(ln[4]) == r["loss"]
