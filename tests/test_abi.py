"""The engine library builds for sm_100a, loads, and exports the C ABI.

No compute is launched here (no GPU needed)."""
import ctypes
import os
import subprocess

from rwig_b200 import _lib


def test_header_declares_entry_points():
    syms = _lib.header_symbols()
    for name in ("rwig_init", "rwig_last_error", "rwig_sinkhorn_log", "rwig_sinkhorn_log_dev"):
        assert name in syms


def test_library_exports_every_header_symbol(engine):
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in _lib.header_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # every typed signature in the binding refers to a declared symbol
    assert set(_lib.SIGNATURES) <= set(_lib.header_symbols())


def test_only_c_abi_is_exported(engine):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert exported == set(_lib.header_symbols()), exported ^ set(_lib.header_symbols())


def test_version_and_error_string_without_device(engine):
    assert engine.rwig_version() == 100
    assert isinstance(engine.rwig_last_error(), bytes)


def test_sm100a_only():
    """The build compiles for sm_100a and nothing else."""
    from rwig_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(_lib.LIB_PATH)
