"""The C-ABI library loads and exports every entry point include/bp_b200.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(bp_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared()
    assert "bp_ax_hex3d" in names and "bp_solver_solve" in names and len(names) > 30


def test_library_exports_every_declared_symbol(bp):
    L = bp.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing
    assert set(bp.EXPORTS) == set(_declared())


def test_library_reports_errors_without_gpu_calls(bp):
    # argument validation happens before any device work
    with pytest.raises(bp.BPError, match="degree"):
        d = bp.AxDesc(5, 0, 0, 1)
        bp._check(bp.lib().bp_ax_hex3d(ctypes.byref(d), 1, 1, 1, 1, 1, 1, 1, 1.0, 1, 1, None))
    assert bp.lib().bp_version().decode().startswith("benchparanumal_b200")


def test_library_is_sm100a_only():
    so = os.path.join(ROOT, "benchparanumal_b200", "libbp_b200.so")
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", so], capture_output=True, text=True)
    assert out.returncode == 0
    assert "sm_100a" in out.stdout


def test_cli_help_and_option_errors(bp):
    # -h prints the usage and succeeds without touching a device
    assert bp.driver_main("BP5", ["-h"]) == 0
    # values outside a setting's allowed list abort (settings.cpp updateVal)
    assert bp.driver_main("BP5", ["-p", "16"]) != 0
    assert bp.driver_main("BP5", ["-p", "4", "-p", "5"]) != 0
    assert bp.driver_main("BK5", ["-m", "OpenMP"]) != 0
    assert bp.driver_main("BP9", []) != 0
