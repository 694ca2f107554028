"""The C ABI from C: tests/c_caller.c is compiled as C99 against
include/ct2b200.h (so the header is valid C, not only C++), linked to the
built library, and run without a GPU (it calls only argument checks, empty
inputs and host bookkeeping)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ct-2_b200")


def test_c_caller(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    if not os.path.exists(os.path.join(LIBDIR, "libct2b200.so")):
        pytest.fail("libct2b200.so is not built")
    exe = str(tmp_path / "c_caller")
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_caller.c"), "-o", exe,
                    "-L", LIBDIR, "-lct2b200", "-Wl,-rpath," + LIBDIR],
                   check=True, capture_output=True, text=True)
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    assert "all checks hold" in run.stdout
