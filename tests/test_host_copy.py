"""The multi-threaded host copy out of pinned staging (host_copy.h) covers
every byte of the destination and nothing past it, for sizes with every
remainder, under concurrent callers.  Built with g++ here; no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_copy_covers_every_byte(tmp_path):
    exe = tmp_path / "host_copy_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "jianhui-lbm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "host_copy_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
