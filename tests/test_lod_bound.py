"""The LOD-test certificate of the descent (voxviz_b200/csrc/lod_bound.h):
every level it clears must continue under the exact binary32 test, on random
inputs and on inputs whose pixel size sits one ulp above the exact
projection.  The kernels skip the exact evaluation only at cleared levels,
so their decisions (and the bit-exact parity) rest on this."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_certificate_never_clears_a_stopping_level(tmp_path):
    exe = tmp_path / "lod_bound_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", str(ROOT / "tests" / "lod_bound_check.cpp"),
                    "-o", str(exe)], check=True)
    total = 0
    for seed in (1, 2, 3):
        r = subprocess.run([str(exe), "200000", str(seed)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        checks, violations = map(int, r.stdout.split())
        assert violations == 0
        total += checks
    assert total > 300000, total  # the certificate does clear levels
