"""Host sanitizers (compute-sanitizer is not used on the GPU pool): the CPU
oracle and the host builder of the cubed-sphere tables, compiled with
AddressSanitizer and UndefinedBehaviorSanitizer, run small cases of every
configuration the path supports; the table driver also checks every ghost
and edge entry against the bounds of the arrays the kernels index with it
(tests/sanitize/)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = ["-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
       "-fno-sanitize-recover=undefined", "-ffp-contract=off"]

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")


def _build_and_run(tmp_path, name, sources, extra=()):
    exe = str(tmp_path / name)
    r = subprocess.run(["g++", *SAN, *extra, *[os.path.join(ROOT, s) for s in sources], "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr[-4000:])
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-4000:]
    return r.stdout


def test_tables_in_bounds_under_sanitizers(tmp_path):
    out = _build_and_run(tmp_path, "tables", ["tests/sanitize/tables_driver.cpp",
                                              "exocubed_b200/csrc/geometry.cpp"])
    assert "tables: ok" in out


def test_oracle_under_sanitizers(tmp_path):
    out = _build_and_run(tmp_path, "oracle", ["oracle/exo_oracle.cpp",
                                              "tests/sanitize/oracle_driver.cpp"])
    assert "oracle: ok" in out


def test_fastdiv_exact_under_sanitizers(tmp_path):
    out = _build_and_run(tmp_path, "fastdiv", ["tests/sanitize/fastdiv_driver.cpp"])
    assert "fastdiv: ok" in out
