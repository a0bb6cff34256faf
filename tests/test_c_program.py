"""The C ABI from C: tests/c/bulk_fluid.c, a plain C program that includes
only include/rmpcd.h and links librmpcd_b200.so, builds with gcc (CPU) and
runs a bulk fluid through the entry points a C or Fortran caller uses (GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def build(tmp_path) -> Path:
    import rmpcdmd_b200 as rm

    lib = Path(rm._capi.LIB_PATH)
    exe = tmp_path / "bulk_fluid"
    cmd = [shutil.which("gcc") or "gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", str(ROOT / "include"), str(ROOT / "tests" / "c" / "bulk_fluid.c"), "-o", str(exe),
           "-L", str(lib.parent), "-lrmpcd_b200", f"-Wl,-rpath,{lib.parent}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_program_builds_against_the_header(tmp_path):
    assert build(tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["64", "32"])
def test_c_program_runs(tmp_path, precision):
    exe = build(tmp_path)
    r = subprocess.run([str(exe), precision], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok" in r.stdout
