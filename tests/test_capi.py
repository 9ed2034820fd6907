"""The C-ABI library loads on a machine without a GPU and exports every
function include/echo_gpu.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from echo_gpu import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "echo_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(echo_gpu_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "echo_gpu_init" in names and "echo_gpu_evolve_main" in names
    assert len(names) >= 20


@pytest.mark.parametrize("exact", [False, True])
def test_library_exports_every_symbol(exact):
    path = L.library_path(exact)
    if not os.path.exists(path):
        pytest.skip("library not built")
    lib = ctypes.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) <= set(L.FUNCTIONS), set(declared()) - set(L.FUNCTIONS)


def test_params_struct_layout_matches_c():
    # the ctypes mirror must have the C layout: ibc is int[16][2][3]
    from echo_gpu.params import EchoParams

    p = EchoParams()
    assert ctypes.sizeof(p.ibc) == 16 * 2 * 3 * 4
    assert EchoParams.cfl.offset % 8 == 0
