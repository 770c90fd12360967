"""The C ABI from C itself: include/edp.h compiles as strict C99, and a C
program links libedp_b200 and calls its device-free entry points (ABI
version, status strings), as a cgo or other FFI caller would."""

import subprocess

import pytest
from conftest import ROOT

LIBDIR = ROOT / "exact-depth-peeling_b200/peel_b200"


def test_header_is_c99(tmp_path):
    source = tmp_path / "header.c"
    source.write_text('#include "edp.h"\nint main(void) { return 0; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I", str(ROOT / "include"), "-fsyntax-only", str(source)], check=True)


def test_c_program_links_and_calls(tmp_path):
    if not (LIBDIR / "libedp_b200.so").exists():
        pytest.skip("libedp_b200.so is not built")
    exe = tmp_path / "c_caller"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests/native/c_caller.c"), "-L", str(LIBDIR), "-ledp_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    done = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert done.returncode == 0, done.stderr
    assert done.stdout.split() == ["abi", "5", "metrics", "24", "status", "16"]
