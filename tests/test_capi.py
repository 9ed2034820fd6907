"""The C-ABI library loads on a machine without a GPU and exports every
function include/echo_gpu.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from echo_gpu import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "echo_gpu.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(echo_(?:gpu|batch)_\w+)\s*\(", src)))


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


def test_struct_layouts_match_the_header(tmp_path):
    """Every field offset and struct size of the ctypes mirrors equals what
    a C compiler gives for include/echo_gpu.h."""
    import shutil
    import subprocess

    from echo_gpu import lib as LB
    from echo_gpu.params import EchoParams

    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    structs = {"EchoParams": EchoParams, "EchoEventGrid": LB.EchoEventGrid, "EchoEventStatus": LB.EchoEventStatus,
               "EchoStats": LB.EchoStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for f in cls._fields_:
            lines.append(f'  printf("{name}.{f[0]} %zu\\n", offsetof({name}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == ctypes.sizeof(cls), name
        for f in cls._fields_:
            assert int(got[f"{name}.{f[0]}"]) == getattr(cls, f[0]).offset, (name, f[0])
