"""The C ABI library loads (no GPU needed) and exports every function include/caelix_b200.h
declares; the header compiles as C99."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "caelix_b200.h")
LIB = os.path.join(REPO, "caelix-renderer_b200", "libcaelix_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"CAELIX_API\s+[\w\s\*]+?\b(caelix_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "caelix_light_bvh_build" in names
    assert "caelix_radix_sort_pairs" in names


def test_library_exports_every_declared_function():
    assert os.path.exists(LIB), "libcaelix_b200.so not built (run make -C caelix-renderer_b200)"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_without_gpu():
    import caelix_b200

    v = caelix_b200.library().version()
    assert v.abi == 2


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_header_is_c99(tmp_path):
    src = tmp_path / "abi.c"
    src.write_text('#include "caelix_b200.h"\nint main(void) { CaelixVersion v; caelix_get_version(&v); return 0; }\n')
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), "-c",
                    str(src), "-o", str(tmp_path / "abi.o")], check=True)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_python_structs_match_the_header(tmp_path):
    """Every ctypes struct of the Python mirror has the C header's size and field offsets."""
    import caelix_b200

    structs = [v for k, v in vars(caelix_b200).items()
               if k.startswith("Caelix") and isinstance(v, type) and issubclass(v, ctypes.Structure)]
    assert any(s.__name__ == "CaelixBatchView" for s in structs)
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "caelix_b200.h"', "int main(void) {"]
    for s in structs:
        lines.append(f'printf("{s.__name__} sizeof %zu\\n", sizeof({s.__name__}));')
        for name, _ in s._fields_:
            lines.append(f'printf("{s.__name__} {name} %zu\\n", offsetof({s.__name__}, {name}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            struct, field, value = line.split()
            got[(struct, field)] = int(value)
    for s in structs:
        assert got[(s.__name__, "sizeof")] == ctypes.sizeof(s), s.__name__
        for name, _ in s._fields_:
            assert got[(s.__name__, name)] == getattr(s, name).offset, (s.__name__, name)
