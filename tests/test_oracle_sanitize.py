"""The C restatement (the oracle) built with AddressSanitizer and
UndefinedBehaviorSanitizer and driven through every step path on small grids
by its host harness (oracle/restate/san_main.c): no out-of-bounds access, use
after free, leak or undefined operation.  Runs on the host; no GPU."""
import os
import shutil
import subprocess

import pytest

ORACLE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")


@pytest.mark.skipif(shutil.which("make") is None or shutil.which("gcc") is None, reason="needs make and gcc")
def test_restatement_clean_under_asan_and_ubsan():
    build = subprocess.run(["make", "-C", ORACLE, "sanitize"], capture_output=True, text=True)
    if build.returncode != 0 and "sanitize" in build.stderr and "libasan" in build.stderr:
        pytest.skip("the compiler has no sanitizer runtime")
    assert build.returncode == 0, build.stderr[-2000:]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    run = subprocess.run([os.path.join(ORACLE, "_build", "san", "oracle_san")], capture_output=True, text=True,
                         env=env, timeout=600)
    assert run.returncode == 0, (run.stdout[-2000:], run.stderr[-4000:])
    assert "runtime error" not in run.stderr and "ERROR: AddressSanitizer" not in run.stderr, run.stderr[-4000:]
    assert "0 case(s) failed" in run.stdout
