"""The serving loop's device-pool allocator (adabool_b200/csrc/abf_pool.h),
checked on the host: tests/pool_check.cpp is compiled with g++ and drives it
through random allocations and whole / partial releases against a shadow
list of live ranges."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_pool_allocator_invariants(tmp_path):
    exe = tmp_path / "pool_check"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'adabool_b200' / 'csrc'}",
                    str(ROOT / "tests" / "pool_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
