"""The oracle (and its deck reader) under AddressSanitizer and
UndefinedBehaviorSanitizer: oracle/sanitize_driver.c drives every routine on
a small seeded system from a golden deck; any out-of-bounds access, leak or
undefined behaviour aborts the run."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def test_oracle_clean_under_asan_ubsan(tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("no gcc")
    exe = tmp_path / "sanitize_driver"
    cmd = ["gcc", "-O1", "-g", "-std=c11", "-ffp-contract=off", "-fno-omit-frame-pointer",
           "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           os.path.join(REPO, "oracle", "clmd_oracle.c"),
           os.path.join(REPO, "oracle", "sanitize_driver.c"), "-lm", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([str(exe), os.path.join(HERE, "golden", "nose_vapour.3d")],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "runtime error" not in r.stderr
    assert r.stdout.count("status") == 8
