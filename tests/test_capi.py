"""The C ABI surface: the shared library loads, exports every entry point
the header declares, and the Python mirror keeps the reference's method
names.  No GPU needed."""
import ctypes
import os
import re
import subprocess

import pytest

import mercury_b200 as mb
from mercury_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "mercury_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mb_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = header_functions()
    assert "mb_simulate" in names and "mb_set_elements" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_exports_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mb_\w+)", out))
    assert set(header_functions()) <= exported


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", "-"],
                       input='#include "mercury_b200.h"\nint main(void){return MB_OK;}\n',
                       capture_output=True, text=True, cwd=os.path.join(ROOT, "include"))
    assert r.returncode == 0, r.stderr


def test_version_string():
    assert mb.LIB.mb_version().decode().startswith("mercury_b200")


def test_null_arguments_are_rejected_without_a_device():
    assert mb.LIB.mb_context_create(0, None) == 1  # MB_ERR_ARGUMENT
    assert mb.LIB.mb_set_materials(None, None) == 1
    assert mb.LIB.mb_simulate(None, ctypes.c_float(1.0), 0, None) == 1
    assert mb.LIB.mb_collect(None, None, None, None) == 1
    assert mb.LIB.mb_last_error(None) == b"null context"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_context_without_device_fails_cleanly():
    ctx = ctypes.c_void_p()
    assert mb.LIB.mb_context_create(0, ctypes.byref(ctx)) == 2  # MB_ERR_CUDA, no crash
    assert not ctx.value


def test_python_mirror_keeps_reference_names():
    # class Simulator, Simulator.h:27-48
    for name in ("Initialize", "SetElement", "SetElements", "Simulate", "Devo", "Collect",
                 "CollectElement", "getDeltaT", "setTimeStep", "getTotalTime", "Reset"):
        assert callable(getattr(mb.Simulator, name)), name
    cfg = mb.SimulatorConfig()
    assert (cfg.time_step, cfg.replaced_springs_per_element) == (0.005, 128)  # config.h:16-21


def test_product_does_not_import_the_oracle():
    pkg = os.path.join(ROOT, "mercury_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cpp", ".cu", ".h", ".cuh")):
                src = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in re.sub(r"(#|//).*", "", src).replace("the oracle", ""), f
