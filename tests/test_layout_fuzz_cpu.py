"""The host layout builders under AddressSanitizer and UndefinedBehaviorSanitizer:
20000 random (post, src) tables -- valid, out of range and out of order --
through bt_layout_build and bt_layout_slices (tests/layout_fuzz.cpp checks
every output against a direct construction).  They are the gate of the C
ABI's trust boundary: the device entry points index by what they produce."""

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_layout_builders_under_sanitizers(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    exe = tmp_path / "layout_fuzz"
    build = subprocess.run([cxx, "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined",
                            "-fno-sanitize-recover=all", f"-I{ROOT / 'include'}",
                            str(ROOT / "btorch_b200" / "csrc" / "layout.cpp"), str(ROOT / "tests" / "layout_fuzz.cpp"),
                            "-o", str(exe)], capture_output=True, text=True)
    if build.returncode != 0 and "sanitize" in build.stderr:
        pytest.skip("sanitizer runtime unavailable: " + build.stderr.strip().splitlines()[-1])
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-4000:]
    assert "bad 0" in run.stdout
