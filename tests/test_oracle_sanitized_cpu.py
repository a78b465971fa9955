"""The C oracle itself under AddressSanitizer and UndefinedBehaviorSanitizer:
oracle.c is compiled with both into a temporary library and the golden-vector
tests (tests/test_oracle_golden.py, the reference's own outputs) run again
against it in a child process with the sanitizer runtimes preloaded, so an
out-of-bounds access or undefined operation in the checker fails here instead
of silently corrupting a parity result."""

import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

DRIVER = """
import sys
from pathlib import Path
sys.path.insert(0, {root!r})
import oracle.oracle as O
O.build = lambda force=False: Path({lib!r})
import pytest
sys.exit(pytest.main(["-q", "-x", "-p", "no:cacheprovider", "tests/test_oracle_golden.py"]))
"""


def test_oracle_golden_cases_under_sanitizers(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    runtimes = [subprocess.run([gcc, f"-print-file-name={name}"], capture_output=True, text=True).stdout.strip()
                for name in ("libasan.so", "libubsan.so")]
    if not all(os.path.isabs(r) and os.path.exists(r) for r in runtimes):
        pytest.skip("sanitizer runtimes unavailable")
    lib = tmp_path / "liboracle_sanitized.so"
    subprocess.run([gcc, "-O1", "-g", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread",
                    "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-o", str(lib),
                    str(ROOT / "oracle" / "oracle.c"), "-lm"], check=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:halt_on_error=1", LD_PRELOAD=":".join(runtimes))
    run = subprocess.run([sys.executable, "-c", DRIVER.format(root=str(ROOT), lib=str(lib))], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=1200)
    assert run.returncode == 0, run.stdout[-3000:] + run.stderr[-3000:]
    assert " passed" in run.stdout
